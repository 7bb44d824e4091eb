"""CPU model of the packed MSV pre-screen (csrc/prescreen.cuh), the checker of
its integer arithmetic: the bound the kernel computes for one (profile,
target) pair, bit for bit.

The pre-screen has no counterpart in the reference (its MSV, src/hmmer/dp.rs:92-145,
is f32 only); what the tests require of it is (1) the kernel computes exactly
this model, and (2) the model's bound is never below the reference's f32 MSV
score, so no pair the reference passes through F1 is dropped.
"""
import ctypes
import math

import numpy as np

Q16 = 512                # cells: units of 2^-9 nat
Q32 = 1 << 20            # specials: units of 2^-20 nat
RHO32 = 8                # 2^-17 nat in units of 2^-20
EFLOOR, EPAD, BEFLOOR = -8192, -16384, -16384
NEG16, NEG32 = -32768, -(1 << 30)
LN2_F32 = np.float32(0.693147182464599609375)

_libm = ctypes.CDLL("libm.so.6")
_libm.logf.restype = ctypes.c_float
_libm.logf.argtypes = [ctypes.c_float]


def quantize(msc, m):
    """Rounded-up int16 scores of columns 1..m (25 rows) and the profile's cap."""
    e = np.asarray(msc, np.float32)[:, 1:m + 1]
    finite = e > np.float32(-1e30)
    u = np.full(e.shape, EFLOOR, np.int64)
    u[finite] = np.maximum(np.ceil((e[finite].astype(np.float64) + 2.0 ** -12) * Q16), EFLOOR).astype(np.int64)
    emax = max(EFLOOR, int(u[finite].max())) if finite.any() else EFLOOR
    return u, 32767 - emax, emax


def _q32_up(x):
    """f32 constant x in units of 2^-20 nat, rounded up, plus rho (the device's q32_up)."""
    return int(math.ceil(float(np.float32(x)) * Q32)) + RHO32


def _f32_round_up(v):
    f = np.float32(v)
    if float(f) < v:
        f = np.nextafter(f, np.float32(np.inf))
    return f


def msv_bound(msc, m, msv_tbm, width, dsq):
    """The pre-screen's bound (f32 nats) for one pair; inf when a row maximum
    exceeded the cap; NaN for an empty target.  `width` = G * C of the
    profile's MSV shape (columns past m are padding with score -32 nats)."""
    L = len(dsq)
    if L == 0:
        return np.float32(np.nan)
    u, cap, emax = quantize(msc, m)
    if emax >= 8192:
        return np.float32(np.nan)
    e = np.full((25, width), EPAD, np.int64)
    e[:, :m] = u
    lf = np.float32(L)
    tloop = _libm.logf(np.float32(lf / (lf + np.float32(3.0))))
    tmove = _libm.logf(np.float32(np.float32(3.0) / (lf + np.float32(3.0))))
    tl, tm = _q32_up(tloop), _q32_up(tmove)
    q_tbm = int(math.ceil((float(np.float32(msv_tbm)) + 2.0 ** -17) * Q32))
    nln2 = int(math.ceil(float(-LN2_F32) * Q32)) + RHO32
    prev = np.full(width, NEG16, np.int64)
    xn, xj = 0, NEG32
    be = max((tm + q_tbm + 2047) >> 11, BEFLOOR)
    for x in dsq:
        shifted = np.empty(width, np.int64)
        shifted[0] = NEG16
        shifted[1:] = prev[:-1]
        cur = e[int(x)] + np.maximum(shifted, be)
        xe = int(cur.max())
        if xe > cap:
            return np.float32(np.inf)
        xj = max(xj + tl, xe * 2048 + nln2)
        xn += tl
        xb = max(xn, xj) + tm
        be = max((xb + q_tbm + 2047) >> 11, BEFLOOR)
        prev = cur
    return np.float32(_f32_round_up(xj + tm) * np.float32(2.0 ** -20))
